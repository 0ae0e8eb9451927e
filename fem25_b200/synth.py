"""Seeded synthetic meshes and models for the fem25 hot path.

The reference reads its mesh from ``<proj>.nodes`` / ``<proj>.mesh``
(``mesh_utils.f:982-1165``, RDMESHBK): per element a domain letter and four
anchor nodes, per anchor node a two-letter class, coordinates, PML depths,
Lame parameters and density.  No public dataset exists for this path, so the
benchmark meshes are generated here with the sizes and value distributions of
the benchmark configurations, seeded with ``numpy.random.Generator(PCG64)``.

Conventions (same as the reference):
  * x to the right, z up, free surface on top (z = 0 before topography).
  * anchor order per element: bottom-left, bottom-right, top-right, top-left
    (counter-clockwise, so the Jacobian is positive, ``cjac.f:115-125``).
  * element domains 'A' (PML), 'E' (Bielak strip), 'I' (interior).
  * anchor classes FL/FR/FB (fixed), FS (free surface), AA/EE/II, BA
    (Bielak/absorbing), BI (Bielak/interior) (``mesh_utils.f:997-1009``).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

TWOPI = 6.2831853071795862


@dataclasses.dataclass
class Mesh:
    nelem: int
    nnpg: int
    nord: int
    ieng: np.ndarray      # int32 [nelem, 4], 1-based
    cdomain: np.ndarray   # uint8 [nelem]
    cnnpg: np.ndarray     # uint8 [nnpg, 2]
    xlocs: np.ndarray
    zlocs: np.ndarray
    xd: np.ndarray
    zd: np.ndarray
    ecoeff: np.ndarray    # float64 [2, nnpg]: lambda row, mu row (ECOEFF(NNPG,2))
    dens: np.ndarray
    xwidth: float
    zwidth: float
    rcoeff: tuple = (1e-4, 1e-4)   # (surface-wave 'S', body-wave 'B'), read_ini.f90:241-250
    dmax: tuple = (0.0, 0.0)
    kappa: tuple = (1.0, 1.0)
    fcent: tuple = (0.0, 0.0)
    nx: int = 0
    nz: int = 0
    # dispersive media (RDMESHBK IDISP > 0, mesh_utils.f:1082-1133): quality
    # factors at the anchors and the reference frequency; 9999 = no damping
    ldisp: bool = False
    qp: np.ndarray | None = None
    qs: np.ndarray | None = None
    freq0: float = 0.0


def dmfrho(vp: np.ndarray) -> np.ndarray:
    """Density (kg/m^3) from Vp (m/s), the reference's own law
    (``gengmask.f90:1418-1447``, DMFRHO)."""
    dcoef = [-21893558144627.e-7, 30290041149786.e-7, -18300316791235.e-7,
             63062641966165.e-8, -13556725156168.e-8, 18616741015779.e-9,
             -15948394116079.e-10, 77924797412933.e-12, -16626306058716.e-13]
    v = np.asarray(vp, dtype=np.float64) / 1000.0
    out = np.empty_like(v)
    hi = v >= 5.93
    mid = (v >= 5.5) & (v < 5.93)
    lo = ~(hi | mid)
    out[hi] = 0.9893 + 0.2891 * v[hi]
    if mid.any():
        p = np.zeros(mid.sum())
        vm = v[mid]
        for ij in range(1, 9):
            p = (p + dcoef[9 - ij]) * vm
        out[mid] = p + dcoef[0]
    out[lo] = 1.7407 * v[lo] ** 0.25
    return out * 1000.0


def gaussian_field(rng, nxa, nza, dx, dz, corr_len):
    """Unit-variance Gaussian random field on the anchor grid with a Gaussian
    correlation of length ``corr_len``, made by FFT-filtering white noise."""
    white = rng.standard_normal((nxa, nza))
    kx = np.fft.fftfreq(nxa, d=dx) * TWOPI
    kz = np.fft.fftfreq(nza, d=dz) * TWOPI
    kk = kx[:, None] ** 2 + kz[None, :] ** 2
    filt = np.exp(-0.25 * kk * corr_len ** 2)
    f = np.real(np.fft.ifft2(np.fft.fft2(white) * filt))
    f -= f.mean()
    sd = f.std()
    return f / sd if sd > 0 else f


def structured_mesh(nx, nz, lx, lz, strip, nord=4, seed=0, jitter=0.0, topo_amp=0.0,
                    topo_wavelength=2000.0):
    """Structured nx x nz quad mesh of [0,lx] x [-lz,0].

    ``strip`` elements on the left, right and bottom form the absorbing
    boundary: the outer ceil(strip/2) are PML ('A'), the inner floor(strip/2)
    the Bielak layer ('E').  ``jitter`` moves interior anchors by a uniform
    fraction of the spacing (rejecting any move that would fold an element),
    ``topo_amp`` adds a sinusoidal surface topography blended linearly with
    depth.  Geometry only; the model is set by ``set_model``."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nxa, nza = nx + 1, nz + 1
    dx, dz = lx / nx, lz / nz
    ix, iz = np.meshgrid(np.arange(nxa), np.arange(nza), indexing="ij")
    x = ix * dx
    z = -lz + iz * dz
    x = x.astype(np.float64)
    z = z.astype(np.float64)
    interior = (ix > 0) & (ix < nx) & (iz > 0) & (iz < nz)
    if jitter > 0.0:
        jx = rng.uniform(-jitter, jitter, size=x.shape) * dx
        jz = rng.uniform(-jitter, jitter, size=z.shape) * dz
        x = np.where(interior, x + jx, x)
        z = np.where(interior, z + jz, z)
    if topo_amp > 0.0:
        phase = rng.uniform(0.0, TWOPI)
        top = topo_amp * np.sin(TWOPI * x[:, -1] / topo_wavelength + phase)
        z = z + top[:, None] * (iz / nz)
    aid = (ix * nza + iz + 1).astype(np.int32)  # anchor id, z fastest

    eix, eiz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    eix = eix.reshape(-1)
    eiz = eiz.reshape(-1)
    ieng = np.stack([aid[eix, eiz], aid[eix + 1, eiz], aid[eix + 1, eiz + 1], aid[eix, eiz + 1]],
                    axis=1).astype(np.int32)
    npml = (strip + 1) // 2
    dist = np.minimum(np.minimum(eix, nx - 1 - eix), eiz)
    dom = np.full(eix.shape, ord("I"), np.uint8)
    dom[dist < strip] = ord("E")
    dom[dist < npml] = ord("A")

    xf = x.reshape(-1)
    zf = z.reshape(-1)
    nnpg = nxa * nza
    # element Jacobian sanity (a folded element would make CJMK_TVI fail)
    if jitter > 0.0 or topo_amp > 0.0:
        xa = xf[ieng - 1]
        za = zf[ieng - 1]
        for xi, eta in ((-1, -1), (1, -1), (1, 1), (-1, 1), (0, 0)):
            dsx = 0.25 * np.array([-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)])
            dse = 0.25 * np.array([-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)])
            j = (xa @ dsx) * (za @ dse) - (xa @ dse) * (za @ dsx)
            if (j <= 0).any():
                raise ValueError("jittered mesh folded an element; lower the jitter")

    # anchor classes
    adom = [set() for _ in range(nnpg)]
    for e in range(ieng.shape[0]):
        for a in ieng[e]:
            adom[a - 1].add(chr(dom[e]))
    cn = np.empty((nnpg, 2), np.uint8)
    ixf = ix.reshape(-1)
    izf = iz.reshape(-1)
    for p in range(nnpg):
        if izf[p] == 0:
            c = "FB"
        elif ixf[p] == 0:
            c = "FL"
        elif ixf[p] == nx:
            c = "FR"
        elif izf[p] == nz:
            c = "FS"
        else:
            s = adom[p]
            if s == {"A"}:
                c = "AA"
            elif s == {"E"}:
                c = "EE"
            elif s == {"I"}:
                c = "II"
            elif "I" in s:
                c = "BI"
            else:
                c = "BA"
        cn[p, 0] = ord(c[0])
        cn[p, 1] = ord(c[1])

    # distance into the PML (anchors)
    xl = npml * dx
    xr = lx - npml * dx
    zb = -lz + npml * dz
    xd = np.maximum(0.0, np.maximum(xl - xf, xf - xr))
    zd = np.maximum(0.0, zb - zf)
    xd[np.abs(xd) < 1e-9] = 0.0
    zd[np.abs(zd) < 1e-9] = 0.0
    mesh = Mesh(nelem=ieng.shape[0], nnpg=nnpg, nord=nord, ieng=np.ascontiguousarray(ieng),
                cdomain=dom, cnnpg=cn, xlocs=xf.copy(), zlocs=zf.copy(), xd=xd, zd=zd,
                ecoeff=np.zeros((2, nnpg)), dens=np.zeros(nnpg), xwidth=float(xd.max()),
                zwidth=float(zd.max()), nx=nx, nz=nz)
    return mesh


def set_model_from_velocities(mesh: Mesh, vp, vs, rho):
    vp = np.asarray(vp, np.float64)
    vs = np.asarray(vs, np.float64)
    rho = np.asarray(rho, np.float64)
    mu = vs * vs * rho
    lam = vp * vp * rho - 2.0 * mu   # RDMESHBK INPTYP=1, mesh_utils.f:1135-1138
    mesh.ecoeff = np.ascontiguousarray(np.stack([lam, mu]))
    mesh.dens = np.ascontiguousarray(rho)


def halfspace_model(mesh: Mesh, seed, vp0=3000.0, vs0=1730.0, rho0=2500.0, sigma=0.02,
                    corr_len=1000.0):
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    nxa, nza = mesh.nx + 1, mesh.nz + 1
    dx = (mesh.xlocs.max() - mesh.xlocs.min()) / mesh.nx
    dz = (mesh.zlocs.max() - mesh.zlocs.min()) / mesh.nz
    g = [gaussian_field(rng, nxa, nza, dx, dz, corr_len).reshape(-1) for _ in range(3)]
    set_model_from_velocities(mesh, vp0 * (1 + sigma * g[0]), vs0 * (1 + sigma * g[1]),
                              rho0 * (1 + sigma * g[2]))


def layered_model(mesh: Mesh, seed, vs_layers=(1200.0, 2500.0, 3500.0), vpvs=1.73, pert=0.05):
    rng = np.random.Generator(np.random.PCG64(seed + 11))
    ztop = 0.0
    zbot = float(mesh.zlocs.min())
    depth = (ztop - mesh.zlocs) / (ztop - zbot)       # 0 at top, 1 at bottom
    layer = np.clip((depth * len(vs_layers)).astype(int), 0, len(vs_layers) - 1)
    vs = np.asarray(vs_layers)[layer]
    vs = vs * (1.0 + pert * rng.uniform(-1.0, 1.0, size=vs.shape))
    vp = vpvs * vs * (1.0 + pert * rng.uniform(-1.0, 1.0, size=vs.shape))
    rho = dmfrho(vp)
    set_model_from_velocities(mesh, vp, vs, rho)


def ky_list(freq, nky, vs_min):
    """nky wavenumbers uniformly spaced on [0, 1.2 omega / Vs_min] mapped to
    apparent slowness py = ky/omega (the operator takes py, estiff25.f:61)."""
    omega = TWOPI * freq
    ky = np.linspace(0.0, 1.2 * omega / vs_min, nky)
    return ky / omega


def vs_min(mesh: Mesh):
    return float(np.sqrt(mesh.ecoeff[1] / mesh.dens).min())


CONFIGS = {
    # plain method, small: 40x20, 20 km x 10 km, 0.5 Hz x 16 ky, strip 2
    0: dict(nx=40, nz=20, lx=20000.0, lz=10000.0, strip=2, model="halfspace",
            freqs=[0.5], nky=[16], nsrc=1, jitter=0.0, topo=0.0),
    # batched assembly: 400x120, 8 f over 0.2-1.6 Hz x 64 ky
    1: dict(nx=400, nz=120, lx=200000.0, lz=60000.0, strip=2, model="layered",
            freqs=list(np.linspace(0.2, 1.6, 8)), nky=[64] * 8, nsrc=0, jitter=0.0, topo=0.0),
    # adjoint gradient: the 400x120 layered mesh, 32 sources, 8 f x 64 ky
    2: dict(nx=400, nz=120, lx=200000.0, lz=60000.0, strip=2, model="layered",
            freqs=list(np.linspace(0.2, 1.6, 8)), nky=[64] * 8, nsrc=32, jitter=0.0, topo=0.0),
    # split-precision contraction: 300x150 jittered, 128 src x 96 ky x 12 f
    3: dict(nx=300, nz=150, lx=150000.0, lz=75000.0, strip=2, model="layered",
            freqs=list(np.linspace(0.2, 2.4, 12)), nky=[96] * 12, nsrc=128, jitter=0.2, topo=0.0),
    # uneven batch: 600x200 jittered, strip 4, topography, 24 f, nky=ceil(16 f/0.1)
    4: dict(nx=600, nz=200, lx=300000.0, lz=100000.0, strip=4, model="layered",
            freqs=[0.1 * (i + 1) for i in range(24)],
            nky=[int(math.ceil(16 * 0.1 * (i + 1) / 0.1 - 1e-9)) for i in range(24)],
            nsrc=64, jitter=0.2, topo=200.0),
}


def make_dispersive(mesh: Mesh, seed: int, freq0: float = 1.0, qs_mean: float = 40.0) -> Mesh:
    """Turn ``mesh`` into a dispersive medium: Qs around ``qs_mean`` with a
    seeded +-25 % variation, Qp = 2.25 Qs (the common Qp/Qs ratio for a
    Poisson solid), reference frequency ``freq0``; a few anchors keep the
    reference's "no damping" value 9999."""
    rng = np.random.default_rng(seed)
    qs = qs_mean * (1.0 + 0.25 * rng.uniform(-1.0, 1.0, mesh.nnpg))
    qp = 2.25 * qs
    off = rng.random(mesh.nnpg) < 0.05
    qs[off] = 9999.0
    qp[off] = 9999.0
    mesh.qp, mesh.qs, mesh.freq0, mesh.ldisp = qp, qs, float(freq0), True
    return mesh


def write_mesh(mesh: Mesh, projnm: str, inptyp: int = 2, latlon=(0.0, 0.0, 0.0, 1.0)) -> None:
    """Writes PROJNM.nodes and PROJNM.mesh in the layout RDMESHBK reads
    (``mesh_utils.f:982-1165``): element records (CDOMAIN, IENG(1:4)), then a
    header (NNPG, INPTYP, NORD, IITYPE=1, IDISP), the Bielak/absorbing corner
    coordinates and anchor records (CNNPG, X, Z, XD, ZD, model, DENS [, QP,
    QS]).  inptyp 2 writes (lambda, mu) exactly (shortest round-trip decimal);
    inptyp 1 writes (Vp, Vs)."""
    with open(projnm + ".nodes", "w") as f:
        f.write(f"{mesh.nelem}\n")
        for e in range(mesh.nelem):
            i = mesh.ieng[e]
            f.write(f"'{chr(mesh.cdomain[e])}' {i[0]} {i[1]} {i[2]} {i[3]}\n")
    idisp = 1 if mesh.ldisp else 0
    with open(projnm + ".mesh", "w") as f:
        f.write(f"{mesh.nnpg} {inptyp} {mesh.nord} 1 {idisp}\n")
        f.write(" ".join(repr(float(x)) for x in latlon) + "\n")
        lam, mu, rho = mesh.ecoeff[0], mesh.ecoeff[1], mesh.dens
        for p in range(mesh.nnpg):
            if inptyp == 1:
                model = (np.sqrt((lam[p] + 2.0 * mu[p]) / rho[p]), np.sqrt(mu[p] / rho[p]))
            else:
                model = (lam[p], mu[p])
            vals = [mesh.xlocs[p], mesh.zlocs[p], mesh.xd[p], mesh.zd[p], *model, rho[p]]
            if mesh.ldisp:
                vals += [mesh.qp[p], mesh.qs[p]]
            cls = bytes(mesh.cnnpg[p]).decode()
            f.write(f"'{cls}' " + " ".join(repr(float(v)) for v in vals) + "\n")


def make_config(idx, nx=None, nz=None):
    """Mesh + model + (freq, py) pairs for benchmark configuration ``idx``.
    ``nx``/``nz`` override the element counts (same physical size), for
    small-scale tests of the same configuration."""
    c = CONFIGS[idx]
    nx = c["nx"] if nx is None else nx
    nz = c["nz"] if nz is None else nz
    seed = 2025 + idx
    mesh = structured_mesh(nx, nz, c["lx"], c["lz"], c["strip"], seed=seed,
                           jitter=c["jitter"], topo_amp=c["topo"])
    if c["model"] == "halfspace":
        halfspace_model(mesh, seed)
    else:
        layered_model(mesh, seed)
    vmin = vs_min(mesh)
    pairs = []
    for f, nk in zip(c["freqs"], c["nky"]):
        for py in ky_list(f, nk, vmin):
            pairs.append((float(f), float(py)))
    return mesh, pairs, c


def dof_coords(mesh: Mesh, g) -> tuple[np.ndarray, np.ndarray]:
    """(x, z) of every DOF: the element's GLL node (ILXI, ILETA)
    (node IAE = (ILETA-1) NLXI + ILXI, dshl.f:41-62) mapped through the
    bilinear anchor map (csf2d.f:45-66).  Fixed DOFs (LM = 0) are skipped."""
    nl = mesh.nord + 1
    gll = {4: np.array([-1.0, -math.sqrt(3.0 / 7.0), 0.0, math.sqrt(3.0 / 7.0), 1.0])}.get(
        mesh.nord)
    if gll is None:
        raise ValueError("dof_coords: GLL nodes tabulated for NORD = 4 only")
    xi = np.tile(gll, nl)
    eta = np.repeat(gll, nl)
    sf = 0.25 * np.stack([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta),
                          (1 - xi) * (1 + eta)], axis=1)            # [nen, 4]
    xe = mesh.xlocs[mesh.ieng - 1] @ sf.T                          # [nelem, nen]
    ze = mesh.zlocs[mesh.ieng - 1] @ sf.T
    x = np.zeros(g.ndof)
    z = np.zeros(g.ndof)
    lm = np.asarray(g.lm)                                          # [nelem, nen, 3]
    for c in range(3):
        d = lm[:, :, c].reshape(-1)
        keep = d > 0
        x[d[keep] - 1] = xe.reshape(-1)[keep]
        z[d[keep] - 1] = ze.reshape(-1)[keep]
    return x, z


def smooth_fields(mesh: Mesh, g, pairs, nsrc: int, seed: int, device="cpu", speed=2500.0,
                  corr_len=5000.0, sigma_amp=0.1, nmodes=64):
    """Seeded complex128 nodal fields [len(pairs), nsrc, NDOF] of the adjoint-
    gradient workload: per (pair, source) a lognormal(0, sigma_amp) amplitude
    times exp(i (k0 x + phi)), k0 = omega / speed along x and phi a smooth
    random phase with a Gaussian correlation of length corr_len (a sum of
    nmodes random Fourier modes), scaled to unit RMS.  Built with torch on
    ``device``."""
    import torch
    x, z = dof_coords(mesh, g)
    gen = torch.Generator(device="cpu")
    gen.manual_seed(seed)
    xt = torch.from_numpy(x).to(device)
    zt = torch.from_numpy(z).to(device)
    out = torch.empty((len(pairs), nsrc, g.ndof), dtype=torch.complex128, device=device)
    # modes are summed in chunks of 16 rows ([16, NDOF] per chunk), a handful
    # of launches per source instead of several per mode
    chunk = 16
    for p, (f, _py) in enumerate(pairs):
        k0 = TWOPI * f / speed
        for s in range(nsrc):
            kx = (torch.randn(nmodes, generator=gen, dtype=torch.float64) / corr_len).to(device)
            kz = (torch.randn(nmodes, generator=gen, dtype=torch.float64) / corr_len).to(device)
            b = (torch.rand(nmodes, generator=gen, dtype=torch.float64) * TWOPI).to(device)
            phi = torch.zeros(g.ndof, dtype=torch.float64, device=device)
            for m0 in range(0, nmodes, chunk):
                sl = slice(m0, min(nmodes, m0 + chunk))
                arg = torch.outer(kx[sl], xt)
                arg.addcmul_(kz[sl, None], zt[None, :]).add_(b[sl, None])
                phi += torch.cos_(arg).sum(0)
            phi *= math.sqrt(2.0 / nmodes)
            amp = torch.exp(sigma_amp * torch.randn(g.ndof, generator=gen,
                                                    dtype=torch.float64).to(device))
            v = amp * torch.exp(1j * (k0 * xt + phi))
            out[p, s] = v / torch.sqrt(torch.mean(torch.abs(v) ** 2))
    return out
