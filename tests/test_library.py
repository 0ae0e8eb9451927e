"""CPU checks of the product library: it loads, exports every entry point of
include/fem25gpu.h, and its host-side graph builder (GEN_GRAPH25) is
bit-identical to the oracle's on structured, jittered and topographic meshes."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from fem25_b200 import graph_build, lib, synth

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
