"""CPU checks of the product library: it loads, exports every entry point of
include/fem25gpu.h, and its host-side graph builder (GEN_GRAPH25) is
bit-identical to the oracle's on structured, jittered and topographic meshes."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from fem25_b200 import fazmod, graph_build, lib, read_mesh, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "fem25gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void)\s+(fem25_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_header():
    L = lib()
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
        assert isinstance(getattr(L, s), ctypes._CFuncPtr)


def test_fortran_module_binds_header_symbols():
    """Every BIND(C, NAME=...) of the ISO_C_BINDING module names an entry point
    of the header that the library exports, with the header's argument count."""
    src = open(os.path.join(ROOT, "fortran", "fem25gpu_mod.f90")).read()
    hdr = open(os.path.join(ROOT, "include", "fem25gpu.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    binds = re.findall(r"(?:FUNCTION|SUBROUTINE)[ \t]+\w+\(([^)]*)\)[^\n]*(?:\n[^\n]*?)??"
                       r"BIND\(C,\s*NAME='(fem25_\w+)'\)", src)
    assert len(binds) >= 12
    L = lib()
    for args, name in binds:
        assert hasattr(L, name), name
        m = re.search(r"(?:int|void)\s+" + name + r"\s*\(([^)]*)\)", hdr)
        assert m, name
        nargs_c = len([a for a in m.group(1).split(",") if a.strip()])
        nargs_f = len([a for a in args.replace("&", " ").split(",") if a.strip()])
        assert nargs_c == nargs_f, (name, nargs_c, nargs_f)


@pytest.mark.parametrize("idx,kw", [(0, {}), (1, dict(nx=24, nz=8)), (3, dict(nx=20, nz=10)),
                                    (4, dict(nx=30, nz=12))])
def test_graph_matches_oracle(idx, kw):
    mesh, _, _ = synth.make_config(idx, **kw)
    go = oracle.graph_build(mesh)
    gp = graph_build(mesh)
    assert (go.nnp, go.ndof, go.nzero) == (gp.nnp, gp.ndof, gp.nzero)
    for k in ("ien", "lm", "irptr", "jcptr", "cnp"):
        assert np.array_equal(getattr(go, k), getattr(gp, k)), k


def test_graph_rejects_bad_mesh():
    mesh, _, _ = synth.make_config(0, nx=6, nz=4)
    mesh.ieng = mesh.ieng.copy()
    mesh.ieng[3, 1] = mesh.nnpg + 5
    with pytest.raises(Exception):
        graph_build(mesh)


def test_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from fem25_b200 import Context, Fem25Error
    mesh, _, _ = synth.make_config(0, nx=6, nz=4)
    with pytest.raises(Fem25Error):
        Context(mesh)


@pytest.mark.parametrize("disp", [False, True])
def test_mesh_files_round_trip(tmp_path, disp):
    """synth.write_mesh -> fem25_read_mesh (RDMESHBK) returns the same arrays
    bit for bit with INPTYP 2, and the graph built from the read mesh equals
    the original's."""
    mesh, _, _ = synth.make_config(4, nx=14, nz=6)
    if disp:
        mesh = synth.make_dispersive(mesh, 5)
    proj = str(tmp_path / "model")
    synth.write_mesh(mesh, proj, latlon=(40.1, -120.5, 40.3, -119.9))
    got, info = read_mesh(proj)
    for k in ("ieng", "cdomain", "cnnpg", "xlocs", "zlocs", "xd", "zd", "ecoeff", "dens"):
        assert np.array_equal(getattr(got, k), getattr(mesh, k)), k
    assert got.xwidth == mesh.xd.max() and got.zwidth == mesh.zd.max()
    assert info["neleme"] == int(np.sum(mesh.cdomain == ord("E")))
    assert info["nabs"] == int(np.sum(mesh.cdomain == ord("A")))
    assert (info["xlatmin"], info["xlonmax"]) == (40.1, -119.9)
    assert got.ldisp == disp
    if disp:
        assert np.array_equal(got.qp, mesh.qp) and np.array_equal(got.qs, mesh.qs)
    g0, g1 = graph_build(mesh), graph_build(got)
    for k in ("ien", "lm", "irptr", "jcptr", "cnp"):
        assert np.array_equal(getattr(g0, k), getattr(g1, k)), k


def test_mesh_files_velocity_input_and_errors(tmp_path):
    """INPTYP 1 (Vp, Vs) becomes mu = Vs^2 rho, lambda = Vp^2 rho - 2 mu;
    missing or truncated files are errors, not crashes."""
    mesh, _, _ = synth.make_config(0, nx=6, nz=4)
    proj = str(tmp_path / "vel")
    synth.write_mesh(mesh, proj, inptyp=1)
    got, info = read_mesh(proj)
    assert info["inptyp"] == 1
    assert np.allclose(got.ecoeff, mesh.ecoeff, rtol=1e-12, atol=0)
    with pytest.raises(Exception):
        read_mesh(str(tmp_path / "missing"))
    lines = open(proj + ".mesh").read().splitlines()
    open(proj + ".mesh", "w").write("\n".join(lines[:-3]) + "\n")
    with pytest.raises(Exception):
        read_mesh(proj)


def test_graph_cache(tmp_path):
    """graph_build(cache=...) writes the graph once, reads it back for the same
    mesh and rebuilds it for another mesh or a corrupt file."""
    mesh, _, _ = synth.make_config(0, nx=8, nz=5)
    path = str(tmp_path / "g.bin")
    g0 = graph_build(mesh, cache=path)
    assert os.path.exists(path)
    g1 = graph_build(mesh, cache=path)
    for k in ("ien", "lm", "irptr", "jcptr", "cnp"):
        assert np.array_equal(getattr(g0, k), getattr(g1, k)), k
    other, _, _ = synth.make_config(0, nx=9, nz=5)
    h = ctypes.c_void_p()
    from fem25_b200.lib import _MeshKeep
    mk = _MeshKeep(other)
    assert lib().fem25_graph_load(mk.ptr, os.fsencode(path), ctypes.byref(h)) != 0
    g2 = graph_build(other, cache=str(tmp_path / "g2.bin"))
    assert g2.ndof != g0.ndof
    data = open(path, "rb").read()
    open(path, "wb").write(data[:len(data) // 2])
    mk0 = _MeshKeep(mesh)
    assert lib().fem25_graph_load(mk0.ptr, os.fsencode(path), ctypes.byref(h)) != 0


def test_fazmod_vincenty_published_case():
    """FAZMOD's Vincenty inverse on the published Flinders Peak -> Buninyong
    example (WGS-84 forward azimuth 306 deg 52' 05.37"), plus the same-point
    and due-east / due-north cases."""
    dms = lambda d, m, s: np.sign(d) * (abs(d) + m / 60.0 + s / 3600.0)
    az = fazmod(dms(-37, 57, 3.72030), dms(144, 25, 29.52440), dms(-37, 39, 10.15610),
                dms(143, 55, 35.38390))
    assert abs(az - dms(306, 52, 5.37)) <= 5e-6, az
    assert fazmod(10.0, 20.0, 10.0, 20.0) == 0.0
    assert abs(fazmod(0.0, 0.0, 0.0, 1.0) - 90.0) <= 1e-9
    assert abs(fazmod(0.0, 0.0, 1.0, 0.0) - 0.0) <= 1e-9
